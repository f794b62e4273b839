// Inline-PTX wrappers shared by the kernels that stage data through shared
// memory with mbarriers (sm_100a): barrier set-up, bounded waits, arrivals,
// and 1-D bulk copies from global to shared memory (this GPU's memory only,
// no cluster multicast).
#pragma once

#include <cstdint>

namespace dfb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One poll: true when the phase with the given parity has completed.
__device__ __forceinline__ bool mbar_test(uint64_t* m, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(smem_u32(m)), "r"(parity)
      : "memory");
  return done != 0;
}

// Wait until the phase with the given parity has completed; false after
// `limit` unsuccessful polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* m, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; i++)
    if (mbar_test(m, parity)) return true;
  return false;
}

// The same, giving up early once *stop is set (by a thread that timed out).
__device__ __forceinline__ bool mbar_wait_or_stop(uint64_t* m, uint32_t parity, uint32_t limit,
                                                  const volatile int* stop) {
  for (uint32_t i = 0; i < limit; i++) {
    if (mbar_test(m, parity)) return true;
    if ((i & 63) == 63 && *stop) return false;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* m) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(m)) : "memory");
}

// Arrive and add `bytes` to the transactions the current phase waits for.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* m, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes)
               : "memory");
}

// Bulk copy of `bytes` (a multiple of 16) from global address src (16-byte
// aligned) to shared memory dst (16-byte aligned), completing on mbarrier m.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* m) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(m))
      : "memory");
}

}  // namespace dfb
