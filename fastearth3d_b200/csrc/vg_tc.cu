// Split-precision tensor-core stages of the 3-D viscosity advance (sm_100a).
//
// The pseudo-spectral stress product of advance_memory_3d
// (src/vilma_response.f90:1171-1319, transforms of src/vilma_tensor_sh.f90:168-387)
// is four dense contractions per FE sub-step, each run here on the 5th-generation
// tensor cores (tcgen05.mma kind::tf32, FP32 accumulators in tensor memory) with
// every operand split into two TF32 terms, x = hi + lo, and three products per
// k-step (hi.hi + hi.lo + lo.hi; the dropped lo.lo term is ~2^-22 |a||b|):
//
//   synth    per (order m, product p): S[j][n] = sum_l T_p(l,m; j) X[l][n]
//            equatorial parity halves the work: E (l+m even) and O (l+m odd) sums
//            on the northern rows j < nh, S_j = E + O, S_mirror = sigma_T (E - O)
//   inverse  per latitude j: the longitude inverse DFT of every (p, field) row,
//            split by the half period (phi + pi flips odd m): ev_i (even m >= 2),
//            od_i (odd m) for i = 1..half-1 on the tensor cores, the m = 0 term
//            and the i = 0 column on CUDA cores in FP64; epilogue: times
//            -M(theta_j, phi) dt of the row's element, stored as the even/odd
//            combinations s_i = g_i + g_{i+half}, d_i = g_i - g_{i+half}
//   forward  per latitude j: the forward DFT, even m >= 2 from s, odd m from d,
//            m = 0 on CUDA cores; epilogue applies the analysis-input scales
//   analysis per (m, p): the quadrature adjoints, parity-split like synth
//
// Every CTA computes one 128-row tile against two sub-GEMMs (E/O or even/odd),
// each N <= 128 wide, accumulating into 2 x 128 TMEM columns. Operands are
// staged through shared memory in the canonical no-swizzle K-major layout
// (16-byte core-matrix rows): A (the data) is loaded from HBM two chunks
// ahead into registers and split into hi/lo on the fly; B (Legendre tables
// and DFT twiddles) is constant and kept pre-split in HBM in exactly the
// shared-memory image, copied per chunk by two TMA bulk copies (cp.async.bulk
// completing on an mbarrier). One elected thread issues the MMAs;
// tcgen05.commit arrives on a per-stage mbarrier that releases the stage
// buffer. The inverse stage's epilogue stages its latitude's viscosity rates
// in the (then idle) stage ring. All waits are bounded by the global timer and
// raise a status bit instead of hanging.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "vg_device.cuh"
#include "vg_internal.cuh"
#include "vg_tcgen05.cuh"

namespace vg {
namespace tc {

constexpr int TM = 128;           // tile rows (MMA M)
constexpr int TN = 128;           // max columns of one sub-GEMM (MMA N)
constexpr int KC = 16;            // K per pipeline chunk = two tf32 k-steps
constexpr int NSTAGE = 3;         // shared-memory ring depth
constexpr int NTHR = 256;             // loader threads (A operand: fetch, split, store)
constexpr int MMA_WARP = NTHR / 32;   // the warp after them issues the MMAs
constexpr int NTHR_ALL = NTHR + 32;
constexpr int A_WORDS = TM * KC;  // one split term of the A chunk (32-bit words)
constexpr int B_WORDS = TN * KC;
constexpr int STAGE_WORDS = 2 * A_WORDS + 2 * B_WORDS;
constexpr int TMEM_COLS = 256;
constexpr int MAX_L = 511;  // synthesis slot table in shared memory: lmax + 1 entries
constexpr size_t SMEM_BYTES = (size_t)NSTAGE * STAGE_WORDS * 4 + 1024 + 256 + 4 * TM * 8 + (MAX_L + 1) * 4;
constexpr unsigned long long WAIT_NS = 2000000000ull;  // 2 s bound on any wait

enum { ST_SYNTH = 0, ST_INV = 1, ST_FWD = 2, ST_ANA = 3 };

// pre-split operand image of one (batch key, sub-GEMM, N tile)
struct ImgInfo {
  long long off;  // float offset of the hi image; lo follows after kpad * npad words
  int kpad, npad, nvalid, kvalid;
};

struct Args {
  int L, nlat, nh, nphi, half, F, NC, NCOL, nk, ne3d;
  int nts, nti, ntf, nta;  // N tiles per stage
  const int* kbeg;
  const float* X;     // [(nk + 1)][4][NC]
  float* S;           // [M][nlat][6][NC]   synthesis products, later the analysis inputs
  float* Gs;          // [nlat][2][half][NCOL]
  float* dy;          // [(nk + 1)][6][NC]
  const float* rate;  // [nlat][nphi][ne3d]  mu / eta_eff
  float dt;
  int trap;  // trapezoidal scheme: the factor M / (1 + M/2) instead of M
  const double* invsin;
  const float* img;
  const ImgInfo* info;
  unsigned long long* status;
};

// ------------------------------------------------------------------ PTX helpers
// (shared ones in vg_tcgen05.cuh)
using namespace vg::ptx;

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// bounded waits of this file: the fixed 2 s bound
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity) { return mbar_wait_ns(bar, parity, WAIT_NS); }
__device__ bool mbar_wait_or_abort(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  return mbar_wait_or_abort_ns(bar, parity, abort_flag, WAIT_NS);
}

// instruction descriptor: F32 accumulate, A and B TF32, both K-major
__host__ __device__ constexpr uint32_t idesc_tf32(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
      : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ------------------------------------------------------------------ per-stage geometry

__device__ __forceinline__ int slot_row(const int* kbeg, int l, int m, int nk) {
  return l >= 1 ? __ldg(&kbeg[l]) + m : nk;  // read-only: not ordered behind the epilogue's stores
}

// table sign under theta -> pi - theta (times (-1)^(l+m)): P, G even; dP, H odd
__device__ __forceinline__ float table_sigma(int p) { return (p == 1 || p == 5) ? -1.0f : 1.0f; }
__device__ __forceinline__ int table_of(int p) {
  const int t[6] = {0, 1, 0, 0, 2, 3};
  return t[p];
}

struct Cta {
  int rows;           // valid rows in this tile
  int row0;           // first global row
  int batch_m, p, j;  // stage coordinates
  int nt;
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

// Loader context of one thread: the tile row it stages and that row's
// constant base address (computed once per CTA).
struct RowCtx {
  bool live;
  const float* base;
  int p;
  double is_j;  // 1 / sin(theta_j) for the inverse stage's p = 2 rows
};

template <int STAGE>
__device__ __forceinline__ RowCtx row_ctx(const Args& A, const Cta& c, int r) {
  RowCtx rc;
  const int row = c.row0 + r;
  rc.live = r < c.rows;
  rc.p = 0;
  rc.is_j = 0.0;
  if (STAGE == ST_SYNTH) {
    const int chan = (c.p == 0) ? 0 : (c.p <= 2 ? 1 : (c.p == 3 ? 2 : 3));
    rc.base = A.X + (size_t)chan * A.NC + row;  // + slot * 4 NC
  } else if (STAGE == ST_INV) {
    rc.p = row / A.F;
    const int f = row % A.F;
    rc.base = A.S + ((size_t)c.j * 6 + rc.p) * A.NC + 2 * f;  // + m nlat 6 NC
    rc.is_j = A.invsin[c.j];
  } else if (STAGE == ST_FWD) {
    rc.base = A.Gs + (size_t)c.j * 2 * A.half * A.NCOL + row;  // + (sub half + i) NCOL
  } else {
    rc.base = A.S + (size_t)c.batch_m * A.nlat * 6 * A.NC + (size_t)c.p * A.NC + row;  // + j 6 NC
  }
  if (!rc.live) rc.base = nullptr;
  return rc;
}

// raw values of one quad (four consecutive K of one row; the analysis also
// holds the mirrored latitude's four values)
struct Quad {
  float v[8];
};

// Issue the global loads of one quad (zeros outside the valid K range).
template <int STAGE>
__device__ __forceinline__ void fetch(const Args& A, const Cta& c, const RowCtx& rc, const int* slot_sm, int sub,
                                      int k0, Quad& Q) {
#pragma unroll
  for (int i = 0; i < 8; ++i) Q.v[i] = 0.f;
  if (!rc.live) return;
  if (STAGE == ST_SYNTH) {
    // X[slot(l, m)][chan_p][n], l = m + par + 2 kk
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int dl = sub + 2 * (k0 + q);
      if (c.batch_m + dl <= A.L) Q.v[q] = rc.base[(size_t)slot_sm[dl] * 4 * A.NC];
    }
  } else if (STAGE == ST_INV) {
    // (m, re), (m, im), (m + 2, re), (m + 2, im), m = (sub ? 1 : 2) + 2 (k / 2)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int m = (sub ? 1 : 2) + 2 * ((k0 >> 1) + h);
      if (m <= A.L) {
        const float2 z = *reinterpret_cast<const float2*>(rc.base + (size_t)m * A.nlat * 6 * A.NC);
        Q.v[2 * h] = z.x;
        Q.v[2 * h + 1] = z.y;
      }
    }
  } else if (STAGE == ST_FWD) {
    // s_i (sub 0) or d_i (sub 1), i = k
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = k0 + q;
      if (i < A.half) Q.v[q] = rc.base[((size_t)sub * A.half + i) * A.NCOL];
    }
  } else {
    // analysis: R_j and R_mirror over the northern rows j = k
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = k0 + q, jm = A.nlat - 1 - j;
      if (j < A.nh) {
        Q.v[q] = rc.base[(size_t)j * 6 * A.NC];
        if (jm != j) Q.v[4 + q] = rc.base[(size_t)jm * 6 * A.NC];
      }
    }
  }
}

// The quad's four A values from its raw loads. `sum` accumulates the CUDA-core
// side terms (inverse: column i = 0, sum_m 2 Re z_m; forward: order 0, sum_i s_i).
template <int STAGE>
__device__ __forceinline__ float4 finish(const Cta& c, const RowCtx& rc, int sub, int k0, const Quad& Q,
                                         double& sum) {
  if (STAGE == ST_INV) {
    float v[4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float re = Q.v[2 * h], im = Q.v[2 * h + 1];
      if (rc.p == 2) {  // i (m / sin theta) z
        const int m = (sub ? 1 : 2) + 2 * ((k0 >> 1) + h);
        const float a = (float)((double)m * rc.is_j);
        const float t = re;
        re = -a * im;
        im = a * t;
      } else if (rc.p == 5) {  // i z
        const float t = re;
        re = -im;
        im = t;
      }
      v[2 * h] = re;
      v[2 * h + 1] = im;
      sum += 2.0 * (double)re;
    }
    return make_float4(v[0], v[1], v[2], v[3]);
  }
  if (STAGE == ST_FWD) {
    if (sub == 0) sum += (double)Q.v[0] + (double)Q.v[1] + (double)Q.v[2] + (double)Q.v[3];
    return make_float4(Q.v[0], Q.v[1], Q.v[2], Q.v[3]);
  }
  if (STAGE == ST_ANA) {  // E: R_j + sigma R_mirror; O: R_j - sigma R_mirror
    const float sg = table_sigma(c.p) * (sub ? -1.0f : 1.0f);
    return make_float4(Q.v[0] + sg * Q.v[4], Q.v[1] + sg * Q.v[5], Q.v[2] + sg * Q.v[6], Q.v[3] + sg * Q.v[7]);
  }
  return make_float4(Q.v[0], Q.v[1], Q.v[2], Q.v[3]);
}

__device__ __forceinline__ void store_split(uint32_t* hi_plane, uint32_t* lo_plane, size_t at, float4 v) {
  uint4 hi, lo;
  hi.x = to_tf32(v.x);
  lo.x = to_tf32(v.x - __uint_as_float(hi.x));
  hi.y = to_tf32(v.y);
  lo.y = to_tf32(v.y - __uint_as_float(hi.y));
  hi.z = to_tf32(v.z);
  lo.z = to_tf32(v.z - __uint_as_float(hi.z));
  hi.w = to_tf32(v.w);
  lo.w = to_tf32(v.w - __uint_as_float(hi.w));
  *reinterpret_cast<uint4*>(hi_plane + at) = hi;
  *reinterpret_cast<uint4*>(lo_plane + at) = lo;
}

// ------------------------------------------------------------------ kernel

template <int STAGE>
__global__ void __launch_bounds__(NTHR_ALL, 2) k_tc_stage(Args A) {
  extern __shared__ unsigned char smraw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
  uint32_t* stage_base = (uint32_t*)sm;
  uint64_t* bars = (uint64_t*)(sm + (size_t)NSTAGE * STAGE_WORDS * 4);  // NSTAGE + 1: MMA done per stage, drain
  uint64_t* bfull = bars + NSTAGE + 1;                                      // NSTAGE: B bulk copy landed
  uint64_t* afull = bfull + NSTAGE;                                         // NSTAGE: A stored by all loaders
  uint32_t* tslot = (uint32_t*)(afull + NSTAGE);
  volatile int* abort_flag = (volatile int*)(tslot + 1);
  double* rsum = (double*)(sm + (size_t)NSTAGE * STAGE_WORDS * 4 + 256);  // [2 subs][2 halves][TM]
  int* slot_sm = (int*)(rsum + 4 * TM);                                     // synthesis: slot(m + dl, m)

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const Cta c = cta_info<STAGE>(A);
  if (c.rows <= 0) return;

  if (tid == 0) {
    for (int i = 0; i <= NSTAGE; ++i) mbar_init(&bars[i], 1);
    for (int i = 0; i < NSTAGE; ++i) mbar_init(&bfull[i], 1);
    for (int i = 0; i < NSTAGE; ++i) mbar_init(&afull[i], NTHR);
    fence_mbar_init();
    *abort_flag = 0;
  }
  if (warp == 0) tmem_alloc(tslot, TMEM_COLS);
  for (int i = tid; i < 4 * TM; i += NTHR_ALL) rsum[i] = 0.0;
  if (STAGE == ST_SYNTH)
    for (int dl = tid; dl <= A.L - c.batch_m; dl += NTHR_ALL)
      slot_sm[dl] = slot_row(A.kbeg, c.batch_m + dl, c.batch_m, A.nk);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  const int nch0 = c.sub[0].kpad / KC, nch1 = c.sub[1].kpad / KC, nch = nch0 + nch1;
  // loader mapping: thread serves row r = tid % TM, quads q = tid / TM + 2 * qq
  const int lr = tid % TM, lh = tid / TM;
  const RowCtx rc = row_ctx<STAGE>(A, c, lr);
  double sum0 = 0.0, sum1 = 0.0;  // loader side sums of the two sub-GEMMs
  constexpr int QPT = (TM * KC / 4) / NTHR;  // quads per thread per chunk
  Quad cur[QPT], nxt[QPT], nx2[QPT];  // A raw loads of chunks ch, ch + 1, ch + 2 (two chunks in flight)
  // B chunk of image `I` (chunk kc) into stage buffer `b`: its hi and lo planes
  // are contiguous runs of npad * KC words in the image (offsets multiples of
  // 64 words), two TMA bulk copies issued by one thread onto bfull[b]
  int b_issued = 0;  // B copies issued (loader thread 0 issues them)
  auto copy_b = [&](int b, const ImgInfo& I, int kc) {
    if (tid == 0) {
      uint32_t* Bhi = stage_base + (size_t)b * STAGE_WORDS + 2 * A_WORDS;
      uint32_t* Blo = Bhi + B_WORDS;
      const uint32_t bytes = (uint32_t)(I.npad * KC * 4);
      const float* src_hi = A.img + I.off + (size_t)kc * KC * I.npad;
      const float* src_lo = src_hi + (size_t)I.kpad * I.npad;
      mbar_expect_tx(&bfull[b], 2 * bytes);
      bulk_g2s(Bhi, src_hi, bytes, &bfull[b]);
      bulk_g2s(Blo, src_lo, bytes, &bfull[b]);
    }
    ++b_issued;
  };
  auto fetch_chunk = [&](int ch, Quad* Q) {
    const int sub = ch < nch0 ? 0 : 1, kc = sub ? ch - nch0 : ch;
#pragma unroll
    for (int qq = 0; qq < QPT; ++qq) fetch<STAGE>(A, c, rc, slot_sm, sub, kc * KC + 4 * (lh + 2 * qq), Q[qq]);
  };
  __shared__ int s_b_issued, s_mma_issued;
  int issued = 0;
  if (warp == MMA_WARP) {
    // ---- MMA issuer: chunk ch once its A (all loaders) and B (bulk copy) landed
    if (lane == 0) {
      int b_done = 0;
      for (int ch = 0; ch < nch; ++ch) {
        const int buf = ch % NSTAGE;
        const uint32_t ph = (uint32_t)((ch / NSTAGE) & 1);
        if (!mbar_wait_or_abort(&afull[buf], ph, abort_flag)) {
          *abort_flag = 1;
          atomicOr(A.status, 1ull << (12 + STAGE));
          break;
        }
        if (!mbar_wait(&bfull[buf], ph)) {
          *abort_flag = 1;
          atomicOr(A.status, 1ull << (4 + STAGE));
          break;
        }
        ++b_done;
        tc_fence_after();
        const int sub = ch < nch0 ? 0 : 1, kc = sub ? ch - nch0 : ch;
        const ImgInfo& I = c.sub[sub];
        uint32_t* Ahi = stage_base + (size_t)buf * STAGE_WORDS;
        uint32_t* Alo = Ahi + A_WORDS;
        uint32_t* Bhi = Alo + A_WORDS;
        uint32_t* Blo = Bhi + B_WORDS;
        const uint32_t idesc = idesc_tf32(TM, I.npad);
        const uint32_t d = tmem + (uint32_t)(sub * TN);
#pragma unroll
        for (int ks = 0; ks < KC / 8; ++ks) {
          const uint32_t aoff = (uint32_t)ks * 2 * TM * 16, boff = (uint32_t)ks * 2 * I.npad * 16;
          const uint64_t dah = sdesc(saddr(Ahi) + aoff, TM * 16, 128);
          const uint64_t dal = sdesc(saddr(Alo) + aoff, TM * 16, 128);
          const uint64_t dbh = sdesc(saddr(Bhi) + boff, I.npad * 16, 128);
          const uint64_t dbl = sdesc(saddr(Blo) + boff, I.npad * 16, 128);
          mma_tf32(d, dah, dbh, idesc, (kc > 0 || ks > 0) ? 1u : 0u);
          mma_tf32(d, dah, dbl, idesc, 1u);
          mma_tf32(d, dal, dbh, idesc, 1u);
        }
        mma_commit(&bars[buf]);
        ++issued;
      }
      if (issued > 0) mma_commit(&bars[NSTAGE]);  // drain: tracks every MMA this thread issued
      s_b_issued = b_done;  // the B copies this side has seen land
      s_mma_issued = issued;
    }
    __syncwarp();
  } else {
    // ---- loaders: A of chunk ch into stage buffer ch % NSTAGE, B bulk copies one chunk ahead
    if (nch > 0) {
      copy_b(0, c.sub[0].kpad > 0 ? c.sub[0] : c.sub[1], 0);
      fetch_chunk(0, cur);
    }
    if (nch > 1) fetch_chunk(1, nxt);
    for (int ch = 0; ch < nch; ++ch) {
      const int buf = ch % NSTAGE;
      const int sub = ch < nch0 ? 0 : 1, kc = sub ? ch - nch0 : ch;
      const bool more = ch + 1 < nch;
      if (more) {
        // stage buffer of chunk ch + 1 was last read by the MMAs of chunk ch + 1 - NSTAGE
        const int nb = (ch + 1) % NSTAGE;
        if (ch + 1 >= NSTAGE && !mbar_wait_or_abort(&bars[nb], (uint32_t)(((ch + 1) / NSTAGE - 1) & 1), abort_flag)) {
          *abort_flag = 1;
          atomicOr(A.status, 1ull << STAGE);
        }
        if (*abort_flag) break;
        const int sub1 = (ch + 1) < nch0 ? 0 : 1, kc1 = sub1 ? ch + 1 - nch0 : ch + 1;
        copy_b(nb, c.sub[sub1], kc1);
      }
      if (ch + 2 < nch) fetch_chunk(ch + 2, nx2);
      // A of chunk ch: finish the loads issued two chunks earlier, split, store
      uint32_t* Ahi = stage_base + (size_t)buf * STAGE_WORDS;
      uint32_t* Alo = Ahi + A_WORDS;
#pragma unroll
      for (int qq = 0; qq < QPT; ++qq) {
        const int q = lh + 2 * qq;
        double part = 0.0;
        const float4 v = finish<STAGE>(c, rc, sub, kc * KC + 4 * q, cur[qq], part);
        if (sub)
          sum1 += part;
        else
          sum0 += part;
        store_split(Ahi, Alo, ((size_t)q * TM + lr) * 4, v);
      }
      fence_async_smem();  // this thread's A stores, visible to the tensor cores
      mbar_arrive(&afull[buf]);
      if (more) {
#pragma unroll
        for (int qq = 0; qq < QPT; ++qq) {
          cur[qq] = nxt[qq];
          nxt[qq] = nx2[qq];
        }
      }
    }
  }
  __syncthreads();
  // B copies still in flight after an abort: wait for them (bounded) before
  // the stage ring is reused or the CTA exits
  if (tid == 0)
    for (int q = s_b_issued; q < b_issued; ++q)
      if (!mbar_wait(&bfull[q % NSTAGE], (uint32_t)((q / NSTAGE) & 1))) atomicOr(A.status, 1ull << (4 + STAGE));
  // drain: the issuer's last commit completes once every MMA has
  bool ok = (*abort_flag == 0);
  if (s_mma_issued > 0 && !mbar_wait(&bars[NSTAGE], 0)) {
    ok = false;
    atomicOr(A.status, 1ull << (8 + STAGE));
  }
  // per-row side sums of the two loader threads
  if (tid < NTHR) {
    rsum[(0 * 2 + lh) * TM + lr] = sum0;
    rsum[(1 * 2 + lh) * TM + lr] = sum1;
  }
  ok = __syncthreads_and(ok) != 0;  // the same epilogue decision in every thread
  tc_fence_after();

  if (ok && !*abort_flag) {  // the MMA warp (chalf 2) finds no columns below and only joins the barriers
    const int quad = warp & 3, chalf = warp >> 2;
    const int r = quad * 32 + lane;  // tile row of this thread
    const int row = c.row0 + r;
    const bool live = r < c.rows;
    const uint32_t tbase = tmem + ((uint32_t)(quad * 32) << 16);
    const bool has0 = nch0 > 0, has1 = nch1 > 0;
    const int ncols = max(has0 ? c.sub[0].npad : 0, has1 ? c.sub[1].npad : 0);
    if (STAGE == ST_SYNTH) {
      const int m = c.batch_m, p = c.p;
      const float sg = table_sigma(p);
      for (int cb = chalf * 64; cb < min(ncols, chalf * 64 + 64); cb += 16) {
        float e[16], o[16];
        if (has0) tmem_ld16(tbase + cb, e); else for (int i = 0; i < 16; ++i) e[i] = 0.f;
        if (has1) tmem_ld16(tbase + TN + cb, o); else for (int i = 0; i < 16; ++i) o[i] = 0.f;
        if (!live) continue;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int j = c.nt * TN + cb + i;
          if (j >= A.nh) break;
          const int jm = A.nlat - 1 - j;
          A.S[(((size_t)m * A.nlat + j) * 6 + p) * A.NC + row] = e[i] + o[i];
          if (jm != j) A.S[(((size_t)m * A.nlat + jm) * 6 + p) * A.NC + row] = sg * (e[i] - o[i]);
        }
      }
    } else if (STAGE == ST_INV) {
      const int p = row / A.F, f = row % A.F, e3 = f / 3;
      float c0 = 0.f;  // m = 0 term (weight 1), the real part of z_0
      if (live && p != 2) {
        const float2 z = *reinterpret_cast<const float2*>(A.S + (((size_t)0 * A.nlat + c.j) * 6 + p) * A.NC + 2 * f);
        c0 = (p == 5) ? -z.y : z.x;
      }
      // the latitude's rates mu / eta (nphi x ne3d floats) staged once in the
      // stage ring, free after the main loop (all MMAs have completed)
      const float* rate_g = A.rate + (size_t)c.j * A.nphi * A.ne3d;
      const float* rate_j = rate_g + e3;
      if (A.nphi * A.ne3d <= NSTAGE * STAGE_WORDS) {  // uniform: fits the ring (always at lmax 128)
        float* rate_s = reinterpret_cast<float*>(stage_base);
        for (int t = tid; t < A.nphi * A.ne3d; t += NTHR_ALL) rate_s[t] = __ldg(&rate_g[t]);
        __syncthreads();
        rate_j = rate_s + e3;
      }
      float* gs = A.Gs + (size_t)c.j * 2 * A.half * A.NCOL + row;
      float* gd = gs + (size_t)A.half * A.NCOL;
      auto emit = [&](int i, float ev, float od) {
        float m1 = rate_j[(size_t)i * A.ne3d] * A.dt, m2 = rate_j[(size_t)(i + A.half) * A.ne3d] * A.dt;
        if (A.trap) {
          m1 = m1 / (1.0f + 0.5f * m1);
          m2 = m2 / (1.0f + 0.5f * m2);
        }
        const float g1 = -m1 * (ev + od), g2 = -m2 * (ev - od);
        gs[(size_t)i * A.NCOL] = g1 + g2;
        gd[(size_t)i * A.NCOL] = g1 - g2;
      };
      if (live && c.nt == 0 && chalf == 0) {
        const double sev = rsum[(0 * 2 + 0) * TM + r] + rsum[(0 * 2 + 1) * TM + r];
        const double sod = rsum[(1 * 2 + 0) * TM + r] + rsum[(1 * 2 + 1) * TM + r];
        emit(0, (float)((double)c0 + sev), (float)sod);
      }
      for (int cb = chalf * 64; cb < min(ncols, chalf * 64 + 64); cb += 16) {
        float e[16], o[16];
        if (has0) tmem_ld16(tbase + cb, e); else for (int i = 0; i < 16; ++i) e[i] = 0.f;
        if (has1) tmem_ld16(tbase + TN + cb, o); else for (int i = 0; i < 16; ++i) o[i] = 0.f;
        if (!live) continue;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int ii = 1 + c.nt * TN + cb + i;
          if (ii >= A.half) break;
          emit(ii, e[i] + c0, o[i]);
        }
      }
    } else if (STAGE == ST_FWD) {
      const int p = row / A.F, f = row % A.F;
      const double isj = A.invsin[c.j];
      const float beta_c = (p == 3 || p == 4) ? 2.0f : (p == 5 ? 4.0f : 1.0f);
      auto out = [&](int m) -> float2* {
        return reinterpret_cast<float2*>(A.S + (((size_t)m * A.nlat + c.j) * 6 + p) * A.NC + 2 * f);
      };
      if (live && c.nt == 0 && chalf == 0) {
        // m = 0: F_0 = (2 pi / nphi) sum_i s_i, real
        const double s0 = rsum[0 * TM + r] + rsum[1 * TM + r];
        const float v = (p == 2) ? 0.f : (float)(beta_c * s0 * (2.0 * PI / (double)A.nphi));
        *out(0) = make_float2(v, 0.f);
      }
      for (int sub = 0; sub < 2; ++sub) {
        if (!(sub ? has1 : has0)) continue;
        const int npad = c.sub[sub].npad, nval = c.sub[sub].nvalid;
        for (int cb = chalf * 64; cb < min(npad, chalf * 64 + 64); cb += 16) {
          float v[16];
          tmem_ld16(tbase + sub * TN + cb, v);
          if (!live) continue;
#pragma unroll
          for (int i = 0; i < 16; i += 2) {
            const int kk = c.nt * TN + cb + i;  // (m, re) column; (m, im) follows
            if (kk >= c.nt * TN + nval) break;
            const int m = (sub ? 1 : 2) + 2 * (kk >> 1);
            const float beta = (p == 2) ? (float)((double)m * isj) : beta_c;
            *out(m) = make_float2(beta * v[i], beta * v[i + 1]);
          }
        }
      }
    } else {
      const int m = c.batch_m, p = c.p;
      for (int sub = 0; sub < 2; ++sub) {
        if (!(sub ? has1 : has0)) continue;
        const int npad = c.sub[sub].npad;
        for (int cb = chalf * 64; cb < min(npad, chalf * 64 + 64); cb += 16) {
          float v[16];
          tmem_ld16(tbase + sub * TN + cb, v);
          if (!live) continue;
#pragma unroll
          for (int i = 0; i < 16; ++i) {
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

// One CTA per image: element (k, n) of the K-major B operand, split into
// tf32 hi/lo and written as [k / 4][npad][4] (hi), then the same for lo.
__global__ void k_tc_images(const ImgJob* __restrict__ jobs, float* __restrict__ img, const double* const* tabs,
                            int L, int nlat, int nh, int nphi, int half) {
  const ImgJob J = jobs[blockIdx.x];
  const int kpad = J.info.kpad, npad = J.info.npad;
  uint32_t* hi = reinterpret_cast<uint32_t*>(img + J.info.off);
  uint32_t* lo = hi + (size_t)kpad * npad;
  const double two_pi = 2.0 * PI;
  for (int t = threadIdx.x; t < kpad * npad; t += blockDim.x) {
    const int n = t % npad, k = t / npad;
    double v = 0.0;
    if (n < J.info.nvalid && k < J.info.kvalid) {
      if (J.kind == 0) {  // B[j][kk] = T(l = m + par + 2 kk, m; j)
        const int j = J.n0 + n, l = J.m + J.par + 2 * k;
        const int lm = J.m * (L + 1) - J.m * (J.m - 1) / 2 + (l - J.m);
        v = tabs[J.table][(size_t)lm * nlat + j];
      } else if (J.kind == 1) {  // B[kk][j] = Tw(l = m + par + 2 kk, m; j)
        const int l = J.m + J.par + 2 * (J.n0 + n), j = k;
        const int lm = J.m * (L + 1) - J.m * (J.m - 1) / 2 + (l - J.m);
        v = tabs[4 + J.table][(size_t)lm * nlat + j];
      } else if (J.kind == 2) {  // B[i][(m, ri)] = 2 cos(m phi_i), -2 sin(m phi_i)
        const int i = 1 + J.n0 + n, m = (J.par ? 1 : 2) + 2 * (k >> 1);
        const int t_ = (int)(((long long)m * i) % nphi);
        const double ang = two_pi * (double)t_ / (double)nphi;
        v = (k & 1) ? -2.0 * sin(ang) : 2.0 * cos(ang);
      } else {  // B[(m, ri)][i] = (2 pi / nphi) (cos(m phi_i), -sin(m phi_i))
        const int kk = J.n0 + n, i = k, m = (J.par ? 1 : 2) + 2 * (kk >> 1);
        const int t_ = (int)(((long long)m * i) % nphi);
        const double ang = two_pi * (double)t_ / (double)nphi, scl = two_pi / (double)nphi;
        v = (kk & 1) ? -scl * sin(ang) : scl * cos(ang);
      }
    }
    const float f = (float)v;
    const uint32_t h = to_tf32(f);
    const uint32_t l_ = to_tf32((float)(v - (double)__uint_as_float(h)));
    const size_t o = ((size_t)(k >> 2) * npad + n) * 4 + (k & 3);
    hi[o] = h;
    lo[o] = l_;
  }
}

}  // namespace tc

// ------------------------------------------------------------------ host

namespace {
int round_up(int x, int m) { return (x + m - 1) / m * m; }
}

struct TcPlan {
  tc::Args a;
  int ntile_rows_nc, ntile_rows_col;
  DArr<float> X, S, Gs, dy, rate, img;
  DArr<tc::ImgInfo> info_synth, info_ana, info_inv, info_fwd;
};

static void tc_release(void* p) { delete static_cast<TcPlan*>(p); }

void visc3d_tc_enable(vg_handle* h) {
  const Grid& G = h->grid;
  cudaStream_t s = h->stream;
  const int L = G.lmax, nlat = G.nlat, nphi = G.nphi, half = nphi / 2;
  if (G.mmax != L) throw Error("vg_enable_visc3d: the tensor-core path needs mmax = lmax");
  if (L > tc::MAX_L) throw Error("vg_enable_visc3d: the tensor-core path supports lmax <= 511");
  const int nh = (nlat + 1) / 2;
  const int F = 3 * h->ne3d, NC = 2 * F, NCOL = 6 * F;
  auto* P = new TcPlan();
  h->tc_plan = P;
  h->tc_plan_release = tc_release;
  tc::Args& a = P->a;
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
  const int TN = tc::TN, KC = tc::KC;
  a.nts = (nh + TN - 1) / TN;
  const int kev = 2 * (L / 2), kod = 2 * ((L + 1) / 2);  // (m, re/im) counts: even m >= 2, odd m
  a.nti = std::max(1, (half - 1 + TN - 1) / TN);
  a.ntf = std::max(1, (std::max(kev, kod) + TN - 1) / TN);
  a.nta = ((L / 2 + 1) + TN - 1) / TN;
  // image jobs
  std::vector<tc::ImgJob> jobs;
  long long off = 0;
  auto add = [&](int kind, int table, int m, int par, int n0, int nvalid, int kvalid) {
    tc::ImgJob J;
    J.kind = kind;
    J.table = table;
    J.m = m;
    J.par = par;
    J.n0 = n0;
    J.info.nvalid = std::max(0, nvalid);
    J.info.kvalid = std::max(0, kvalid);
    if (J.info.nvalid == 0 || J.info.kvalid == 0) {
      J.info.kpad = 0;
      J.info.npad = 16;
      J.info.off = 0;
      return J;
    }
    J.info.npad = round_up(J.info.nvalid, 16);  // M = 128 MMAs take N in steps of 16
    J.info.kpad = round_up(J.info.kvalid, KC);
    J.info.off = off;
    off += 2LL * J.info.kpad * J.info.npad;
    off = (off + 63) / 64 * 64;
    jobs.push_back(J);
    return J;
  };
  std::vector<tc::ImgInfo> isyn, iana, iinv(2 * a.nti), ifwd(2 * a.ntf);
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
  P->info_synth.upload(isyn, s);
  P->info_ana.upload(iana, s);
  P->info_inv.upload(iinv, s);
  P->info_fwd.upload(ifwd, s);
  {
    DArr<tc::ImgJob> d_jobs;
    d_jobs.upload(jobs, s);
    const double* tabs_h[8] = {G.d_plm.p, G.d_dplm.p, h->d_G6.p, h->d_H6.p,
                               h->d_wP.p, h->d_wD.p, h->d_wG.p, h->d_wH.p};
    DArr<const double*> d_tabs;
    d_tabs.alloc(8);
    VG_CUDA(cudaMemcpyAsync(d_tabs.p, tabs_h, sizeof(tabs_h), cudaMemcpyHostToDevice, s));
    tc::k_tc_images<<<(int)jobs.size(), 256, 0, s>>>(d_jobs.p, P->img.p, d_tabs.p, L, nlat, nh, nphi, half);
    VG_CUDA(cudaGetLastError());
    VG_CUDA(cudaStreamSynchronize(s));
  }
  // rates transposed to [j][i][element] (FP32), from the (ne3d, nlat, nphi) FP64 copy
  {
    std::vector<double> r3((size_t)h->ne3d * nlat * nphi);
    VG_CUDA(cudaMemcpyAsync(r3.data(), h->d_MkPerDt3.p, r3.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    VG_CUDA(cudaStreamSynchronize(s));
    std::vector<float> rt(r3.size());
    for (int e = 0; e < h->ne3d; ++e)
      for (int j = 0; j < nlat; ++j)
        for (int i = 0; i < nphi; ++i)
          rt[((size_t)j * nphi + i) * h->ne3d + e] = (float)r3[((size_t)e * nlat + j) * nphi + i];
    P->rate.upload(rt, s);
  }
  P->X.alloc((size_t)(h->nk + 1) * 4 * NC);
  P->S.alloc((size_t)G.M * nlat * 6 * NC);
  P->Gs.alloc((size_t)nlat * 2 * half * NCOL);
  P->dy.alloc((size_t)(h->nk + 1) * 6 * NC);
  a.kbeg = h->d_kbeg.p;
  a.X = P->X.p;
  a.S = P->S.p;
  a.Gs = P->Gs.p;
  a.dy = P->dy.p;
  a.rate = P->rate.p;
  a.invsin = G.d_invsin.p;
  a.img = P->img.p;
  a.status = h->d_maxbits.p + 2;
  P->ntile_rows_nc = (NC + tc::TM - 1) / tc::TM;
  P->ntile_rows_col = (NCOL + tc::TM - 1) / tc::TM;
  static std::atomic<bool> attr{false};  // set once; concurrent handles may race to it
  if (!attr) {
    VG_CUDA(cudaFuncSetAttribute(tc::k_tc_stage<tc::ST_SYNTH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::SMEM_BYTES));
    VG_CUDA(cudaFuncSetAttribute(tc::k_tc_stage<tc::ST_INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::SMEM_BYTES));
    VG_CUDA(cudaFuncSetAttribute(tc::k_tc_stage<tc::ST_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::SMEM_BYTES));
    VG_CUDA(cudaFuncSetAttribute(tc::k_tc_stage<tc::ST_ANA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::SMEM_BYTES));
    attr = true;
  }
  VG_CUDA(cudaStreamSynchronize(s));
}

void visc3d_tc_buffers(vg_handle* h, float** X, float** dy) {
  TcPlan* P = static_cast<TcPlan*>(h->tc_plan);
  *X = P->X.p;
  *dy = P->dy.p;
}

// The four tensor-core stages between the FP32 gather and the scatter.
void visc3d_tc_run(vg_handle* h, double dt, bool trap) {
  TcPlan* P = static_cast<TcPlan*>(h->tc_plan);
  const Grid& G = h->grid;
  cudaStream_t s = h->stream;
  tc::Args a = P->a;
  a.dt = (float)dt;
  a.trap = trap ? 1 : 0;
  auto launch = [&](auto kernel, int phase, const tc::ImgInfo* info, dim3 grid) {
    PhaseScope ps(h, phase);
    a.info = info;
    kernel<<<grid, tc::NTHR_ALL, tc::SMEM_BYTES, s>>>(a);
    ++h->n_launch;
    VG_CUDA(cudaGetLastError());
  };
  launch(tc::k_tc_stage<tc::ST_SYNTH>, VG_PH_V3_SYNTH, P->info_synth.p, dim3(P->ntile_rows_nc, a.nts, G.M * 6));
  launch(tc::k_tc_stage<tc::ST_INV>, VG_PH_V3_LON_INV, P->info_inv.p, dim3(P->ntile_rows_col, a.nti, G.nlat));
  launch(tc::k_tc_stage<tc::ST_FWD>, VG_PH_V3_LON_FWD, P->info_fwd.p, dim3(P->ntile_rows_col, a.ntf, G.nlat));
  launch(tc::k_tc_stage<tc::ST_ANA>, VG_PH_V3_ANALYSIS, P->info_ana.p, dim3(P->ntile_rows_nc, a.nta, G.M * 6));
}

}  // namespace vg
