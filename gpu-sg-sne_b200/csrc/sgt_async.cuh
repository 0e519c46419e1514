// sgt_async.cuh -- mbarrier and bulk-copy (TMA engine) helpers shared by the
// kernels that stage global memory into shared memory asynchronously.
// Every wait is bounded: it gives up after SGT_SPIN_CYCLES clock cycles and
// reports that, so a copy that never completes cannot hang the GPU.
#pragma once
#include <cuda_runtime.h>

constexpr long long SGT_SPIN_CYCLES = 4000000000LL;  // clock cycles before a wait gives up

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
// make an initialised mbarrier visible to the async proxy (bulk copies)
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
// bounded wait for the phase with the given parity; false when it gave up
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  const long long t0 = clock64();
  while (true) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > SGT_SPIN_CYCLES) return false;
  }
}
// global -> shared bulk copy into this CTA's own shared memory, completing
// on an mbarrier (both addresses 16-byte aligned, bytes a multiple of 16)
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void *src, unsigned bytes,
                                         unsigned bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}
