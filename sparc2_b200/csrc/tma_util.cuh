// tma_util.cuh -- shared-memory addresses, mbarriers and 3-D / 4-D TMA
// tile loads (cp.async.bulk.tensor, each into the issuing CTA's own shared
// memory), used by the stage and filter kernels.  Every wait on an
// mbarrier is bounded.
#pragma once

#include "internal.h"

namespace sparc {

// polls of an mbarrier before a wait gives up and raises the error flag
constexpr long long kMbarWaitLimit = 1LL << 26;

__device__ __forceinline__ unsigned sm_addr_t(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init_t(unsigned long long *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sm_addr_t(bar)) : "memory");
}
__device__ __forceinline__ void mbar_tx_t(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm_addr_t(bar)),
               "r"(bytes)
               : "memory");
}
// one 3-D tile of the tensor map at (x, y, z) into shared memory at dst,
// completing on bar.  x times the element size must be a multiple of 16
// bytes; coordinates outside the tensor read zero.
__device__ __forceinline__ void tma3d_t(void *dst, const CUtensorMap *map, int x, int y, int z,
                                        unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(sm_addr_t(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(sm_addr_t(bar))
      : "memory");
}
// the same for a 4-D tile at (x, y, z, w)
__device__ __forceinline__ void tma4d_t(void *dst, const CUtensorMap *map, int x, int y, int z,
                                        int w, unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(sm_addr_t(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(sm_addr_t(bar))
      : "memory");
}
// bounded wait: gives up after kMbarWaitLimit polls and raises the error flag
__device__ __forceinline__ bool mbar_wait_t(unsigned long long *bar, unsigned parity, int *err) {
  for (long long n = 0; n < kMbarWaitLimit; ++n) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(sm_addr_t(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  atomicExch(err, 1);
  return false;
}

}  // namespace sparc
