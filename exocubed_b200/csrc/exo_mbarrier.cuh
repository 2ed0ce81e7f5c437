// exo_mbarrier.cuh -- mbarrier and bulk-copy helpers (inline PTX, sm_90+)
// shared by the kernels: a bulk copy global -> shared memory counted on an
// mbarrier, and a wait on an mbarrier phase that gives up after a bounded
// wall time instead of spinning forever.
#pragma once

#include <cuda_runtime.h>

namespace exo {

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* mb, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(mb)), "r"(count)
               : "memory");
}
// one arrival that also announces the bytes the bulk copy will complete
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* mb, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(mb)),
               "r"(bytes)
               : "memory");
}
// bulk copy global -> this CTA's shared memory, counted on mb (no multicast)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         unsigned long long* mb) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(mb))
      : "memory");
}
// Waits for phase `parity` of mb to complete, giving up once MBAR_WAIT_NS of
// wall time (the %globaltimer clock) have passed: false after a timeout.
constexpr unsigned long long MBAR_WAIT_NS = 100000000ull;  // 0.1 s
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_wait(unsigned long long* mb, unsigned parity) {
  const unsigned a = smem_u32(mb);
  const unsigned long long t0 = global_ns();
  for (;;) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (global_ns() - t0 > MBAR_WAIT_NS) return false;
  }
}

}  // namespace exo
