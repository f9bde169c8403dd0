// Inline-PTX helpers of the hand-written tcgen05 kernels (sm_100a): mbarriers
// with bounded waits, tensor-memory allocation, shared-memory matrix
// descriptors, TMA bulk copies (no tensor map, no multicast), MMA commit and
// tensor-memory loads. Shared by the split TF32 stages (vg_tc.cu) and the
// exact int8 stages (vg_oz.cu) of the 3-D viscosity advance.
#pragma once
#include <cstdint>

namespace vg {
namespace ptx {

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Clock of the wait limits: the SM cycle counter (a register read; the global
// timer is a slower read). A limit of `ns` nanoseconds is 2 ns cycles, at least
// `ns` of wall time at any SM clock up to 2 GHz.
__device__ __forceinline__ long long wclock() { return clock64(); }
__device__ __forceinline__ long long wait_cycles(unsigned long long ns) {
  return (long long)(ns > (1ull << 61) ? (1ull << 62) : 2 * ns);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// one potentially blocking test: the hardware suspends the thread until the
// phase completes or about `hint_ns` have passed (no polling loop, so waiting
// threads take no issue slots and read no timer meanwhile)
__device__ __forceinline__ bool mbar_try_hint(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

constexpr uint32_t WAIT_HINT_NS = 20000;  // one suspended test: at most ~20 us

// bounded wait: false after about wait_ns (the clock is read once per
// suspended test)
__device__ __forceinline__ bool mbar_wait_ns(uint64_t* bar, uint32_t parity, unsigned long long wait_ns) {
  if (mbar_try(bar, parity)) return true;
  const long long t0 = wclock(), lim = wait_cycles(wait_ns);
  while (true) {
    if (mbar_try_hint(bar, parity, WAIT_HINT_NS)) return true;
    if (wclock() - t0 > lim) return false;
  }
}

// bounded wait that also gives up once `abort_flag` is raised (the other side
// of a producer / consumer handoff stopped)
__device__ __forceinline__ bool mbar_wait_or_abort_ns(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                                      unsigned long long wait_ns) {
  if (mbar_try(bar, parity)) return true;
  const long long t0 = wclock(), lim = wait_cycles(wait_ns);
  while (true) {
    if (mbar_try_hint(bar, parity, WAIT_HINT_NS)) return true;
    if (*abort_flag || wclock() - t0 > lim) return false;
  }
}

// the same for waiters that are not on the critical path
__device__ __forceinline__ bool mbar_wait_sleep_ns(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                                   unsigned long long wait_ns) {
  return mbar_wait_or_abort_ns(bar, parity, abort_flag, wait_ns);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(bar)) : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// shared-memory matrix descriptor, canonical K-major layout without swizzle:
// 8-row core matrices of 16-byte rows, SBO between 8-row groups, LBO between
// the two 16-byte K halves of one k-step; version 1 (sm_100)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// TMA bulk copy (no tensor map, no multicast): global -> this CTA's shared
// memory, completing `bytes` on the mbarrier's transaction count
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   saddr(dst)),
               "l"(src), "r"(bytes), "r"(saddr(bar))
               : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
               : "memory");
}

}  // namespace ptx
}  // namespace vg
