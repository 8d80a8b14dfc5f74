// tmem_window.cuh -- tensor memory (TMEM, sm_100a) as per-thread storage
// for the register windows of the stage kernels.
//
// The z derivatives of a column use an 11-deep window of values per field,
// three windows per thread.  In FP64 these 33 values take 66 of the 128
// registers a thread of a 512-thread CTA may hold, for the whole layer
// loop.  Kept in TMEM instead, they occupy registers only while the z
// derivatives are formed: each layer loads a window (tcgen05.ld, one wait
// for its three pieces), forms the derivative and stores only the new
// head value (tcgen05.st) into the slot of the layer it replaces, the
// window being a ring whose rotation the caller tracks.  Measured on the
// 256x256x300 flux tube: the FP64 stage kernels lose their register
// spills and run 4.6 % faster (with the whole window stored back shifted
// each layer); storing the head alone into a ring is another 1.1 %; the
// FP32 kernels, which do not spill, ran 4 % slower with their windows in
// TMEM and keep them in registers.
//
// Layout: the CTA (16 warps) allocates all 512 columns.  Warp w may access
// only the lane quarter w % 4 (lanes 32(w%4) .. +31; lane = the thread's
// position in its warp), and the four warps of a quarter take the column
// slices (w / 4) * 128 .. +127.  A thread's windows start at column 0 of
// its slice: fields 0, 1, 2 at 0, 22, 44, a value of 8 bytes in two
// consecutive 32-bit columns (low word first).  The 32-bit columns are
// paired into FP64 registers inside the asm blocks, so no copy of the
// window is held as 32-bit values.  The loads and stores carry no memory
// clobber (they touch no memory the compiler tracks); tm_wait_st orders a
// store before a later load of the same columns.
//
// Every instruction here is warp-collective (.sync.aligned): callers issue
// them with the whole warp converged.  Allocation: one warp allocates and
// frees; the allocation cannot wait on another CTA because only these
// kernels allocate TMEM and two of their CTAs never share an SM (each uses
// the whole register file and more than half of the shared memory).
#pragma once

#include <cstdint>

namespace sparc {

__device__ __forceinline__ uint32_t tm_smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// all 512 columns to the CTA; the TMEM address is written to *slot
__device__ __forceinline__ void tm_alloc_all(uint32_t *slot) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   tm_smem_u32(slot)),
               "r"(512)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tm_free_all(uint32_t taddr) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(512)
               : "memory");
}

__device__ __forceinline__ void tm_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tm_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tm_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tm_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// this warp's window address: lane quarter w % 4, column slice w / 4
__device__ __forceinline__ uint32_t tm_warp_addr(uint32_t base, int warp) {
  return base + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * 128);
}

// One FP64 window (11 values, 22 columns) of this thread at address ta, in
// pieces of 16, 4 and 2 columns: the three loads, one wait and the pairing
// of the 32-bit columns into FP64 registers in one asm block (the
// registers are valid only after the wait), so a window costs one round
// trip to TMEM.  One window at a time keeps 22 registers live, not the 66
// of all three.
__device__ __forceinline__ void tm_ld_window(uint32_t ta, double (&o)[11]) {
  asm volatile(
      "{\n"
      ".reg .b32 t0, t1, t2, t3, t4, t5, t6, t7, t8, t9, t10, t11, t12, t13, t14, t15;\n"
      ".reg .b32 u0, u1, u2, u3, u4, u5;\n"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {t0, t1, t2, t3, t4, t5, t6, t7, t8, t9, t10, t11, t12, t13, t14, t15}, [%11];\n"
      "tcgen05.ld.sync.aligned.32x32b.x4.b32 {u0, u1, u2, u3}, [%12];\n"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {u4, u5}, [%13];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      "mov.b64 %0, {t0, t1};\n"
      "mov.b64 %1, {t2, t3};\n"
      "mov.b64 %2, {t4, t5};\n"
      "mov.b64 %3, {t6, t7};\n"
      "mov.b64 %4, {t8, t9};\n"
      "mov.b64 %5, {t10, t11};\n"
      "mov.b64 %6, {t12, t13};\n"
      "mov.b64 %7, {t14, t15};\n"
      "mov.b64 %8, {u0, u1};\n"
      "mov.b64 %9, {u2, u3};\n"
      "mov.b64 %10, {u4, u5};\n"
      "}"
      : "=d"(o[0]), "=d"(o[1]), "=d"(o[2]), "=d"(o[3]), "=d"(o[4]), "=d"(o[5]), "=d"(o[6]),
        "=d"(o[7]), "=d"(o[8]), "=d"(o[9]), "=d"(o[10])
      : "r"(ta + 0u), "r"(ta + 16u), "r"(ta + 20u));
}

// One FP64 window to address ta (completion: tm_wait_st)
__device__ __forceinline__ void tm_st_window(uint32_t ta, const double (&v)[11]) {
  asm volatile(
      "{\n"
      ".reg .b32 t0, t1, t2, t3, t4, t5, t6, t7, t8, t9, t10, t11, t12, t13, t14, t15;\n"
      "mov.b64 {t0, t1}, %1;\n"
      "mov.b64 {t2, t3}, %2;\n"
      "mov.b64 {t4, t5}, %3;\n"
      "mov.b64 {t6, t7}, %4;\n"
      "mov.b64 {t8, t9}, %5;\n"
      "mov.b64 {t10, t11}, %6;\n"
      "mov.b64 {t12, t13}, %7;\n"
      "mov.b64 {t14, t15}, %8;\n"
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {t0, t1, t2, t3, t4, t5, t6, t7, t8, t9, t10, t11, t12, t13, t14, t15};\n"
      "}" ::"r"(ta + 0u),
      "d"(v[0]), "d"(v[1]), "d"(v[2]), "d"(v[3]), "d"(v[4]), "d"(v[5]), "d"(v[6]), "d"(v[7]));
  asm volatile(
      "{\n"
      ".reg .b32 t0, t1, t2, t3;\n"
      "mov.b64 {t0, t1}, %1;\n"
      "mov.b64 {t2, t3}, %2;\n"
      "tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {t0, t1, t2, t3};\n"
      "}" ::"r"(ta + 16u),
      "d"(v[8]), "d"(v[9]));
  asm volatile(
      "{\n"
      ".reg .b32 t0, t1;\n"
      "mov.b64 {t0, t1}, %1;\n"
      "tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {t0, t1};\n"
      "}" ::"r"(ta + 20u),
      "d"(v[10]));
}

// One FP64 value to address ta (completion: tm_wait_st)
__device__ __forceinline__ void tm_st_one(uint32_t ta, double v) {
  asm volatile(
      "{\n"
      ".reg .b32 t0, t1;\n"
      "mov.b64 {t0, t1}, %1;\n"
      "tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {t0, t1};\n"
      "}" ::"r"(ta),
      "d"(v));
}

// column offset of window f (0, 1, 2) in a thread's slice
__device__ __forceinline__ uint32_t tm_window(uint32_t ta, int f) { return ta + 22u * f; }

}  // namespace sparc
