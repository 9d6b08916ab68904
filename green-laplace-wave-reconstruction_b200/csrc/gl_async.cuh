// Bulk asynchronous global -> shared copies completed on an mbarrier
// (sm_90+ `cp.async.bulk`, no multicast) and a bounded wait on them.
//
// A copy moves `bytes` contiguous bytes (both addresses 16-byte aligned,
// size a multiple of 16) and signals the mbarrier's transaction count; the
// consumer threads wait on phase parity 0.  Every wait is bounded by a clock
// budget so that a copy that never lands turns into an error status instead
// of a hung block.
#pragma once
#include <stdint.h>

#include "gl_common.cuh"

namespace gl {

GL_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

GL_D void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
  // make the initialised barrier visible to the async (bulk copy) proxy
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also adds `bytes` to the expected transaction count.
GL_D void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

GL_D void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// Completes `bytes` of the expected transaction count without a copy.
GL_D void mbar_complete_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.complete_tx.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

GL_D bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

// Wait for phase `parity` for at most `max_cycles` SM clocks.
GL_D bool mbar_wait_bounded(uint32_t bar, uint32_t parity, long long max_cycles) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > max_cycles) return false;
  }
  return true;
}

// ~2 s at the B200's 1.97 GHz boost clock: far above any copy's latency.
constexpr long long BULK_WAIT_CYCLES = 4000000000LL;

}  // namespace gl
