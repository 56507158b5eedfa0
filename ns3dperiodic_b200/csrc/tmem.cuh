// Tensor memory (TMEM) as per-thread storage: the 32x32b access shape gives
// each thread of a warp one TMEM lane (warp w of a 4-warp CTA owns lanes
// 32 w .. 32 w + 31), so a thread can park 32-bit words in its own lane's
// columns and read them back without touching shared memory.
//
// A CTA allocates its columns once (one warp, tcgen05.alloc), publishes the
// address through shared memory across a CTA barrier, and frees them before
// it exits.  An allocation waits until the SM has free columns.  The CTAs
// that hold columns here wait on nothing else, so they always finish and
// free them; callers also bound the CTAs per SM that can hold columns at
// once so that their columns fit the SM's 512 and no allocation waits.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ns3d {

constexpr uint32_t kTmemColsPerSm = 512;

// warp 0 of the CTA: allocate `ncols` (a power of two, 32..512) and write
// their TMEM address to *dst (shared memory); then give up the right to
// allocate again, so other CTAs on the SM are not held back
__device__ __forceinline__ void tmem_alloc_warp(uint32_t* dst, uint32_t ncols) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// warp 0 of the CTA, after every thread's last TMEM access (and a CTA barrier
// between them, fenced as below)
__device__ __forceinline__ void tmem_dealloc_warp(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// order tcgen05 operations around a CTA barrier
__device__ __forceinline__ void tmem_fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// this thread's 8 words at columns col .. col + 7 of its lane
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(
          taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
      : "memory");
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(taddr)
      : "memory");
}
// the thread's earlier tcgen05.st / tcgen05.ld have completed (loaded
// registers may be read after wait_ld)
__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// TMEM address of lane `lane`, column `col` relative to `base`
__device__ __forceinline__ uint32_t tmem_addr(uint32_t base, int lane, int col) {
  return base + ((uint32_t)lane << 16) + (uint32_t)col;
}

}  // namespace ns3d
