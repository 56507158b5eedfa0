// Bulk tensor copies (TMA) into shared memory, completed on mbarriers.
//
// A copy is described by a tensor map (CUtensorMap, built on the host with
// cuTensorMapEncodeTiled over this GPU's own memory) and issued by one
// thread; its completion is counted in bytes on an mbarrier that the
// consumers wait on.  Every wait here is bounded: after 0.1 s (or kMbarSpins
// failed polls) the waiting thread records an error code and carries on, so a
// broken pipeline ends the kernel with a flagged result instead of a hang.
#pragma once

#include <cuda.h>  // CUtensorMap (types only: the library does not link the driver)
#include <cuda_runtime.h>

#include <cstdint>

namespace ns3d {

// How a bounded wait polls: NS3D_TMA_WAIT 1 with try_wait, which suspends
// the thread until the phase completes or kMbarHintNs have passed (the
// waiting warps then take no issue slots from the warps that compute);
// 0 with the non-blocking test_wait, kMbarFast polls back to back, then
// polls spaced by __nanosleep(kMbarSleepNs).  Either way a wait gives up
// after kMbarLimitNs of the global timer, or after kMbarSpins polls.
#ifndef NS3D_TMA_WAIT
#define NS3D_TMA_WAIT 1
#endif
constexpr int kMbarSpins = 1 << 20;
constexpr int kMbarFast = 1 << 10;
constexpr unsigned kMbarSleepNs = 100;
constexpr unsigned kMbarHintNs = 1000;
constexpr unsigned long long kMbarLimitNs = 100000000ull;  // 0.1 s
constexpr int kErrTimeout = 0x54494d45;  // written to the error flag by a wait that gave up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// makes the initialised barriers visible to the async proxy (the TMA unit)
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// the issuing thread's arrival, announcing `bytes` of copies on this phase
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// true once the barrier's phase with this parity has completed (non-blocking)
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// true once the phase with this parity has completed; may suspend the thread
// for up to hint_ns before it returns false
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Polls until the phase completes (true) or the limits of a bounded wait
// pass (false).
__device__ __forceinline__ bool mbar_poll(uint64_t* bar, uint32_t parity) {
  const unsigned long long t0 = global_ns();
  for (int i = 0; i < kMbarSpins; ++i) {
    if (NS3D_TMA_WAIT) {
      if (mbar_try_wait(bar, parity, kMbarHintNs)) return true;
    } else {
      if (mbar_test_wait(bar, parity)) return true;
      if (i >= kMbarFast) __nanosleep(kMbarSleepNs);
    }
    if ((i & 63) == 63 && global_ns() - t0 > kMbarLimitNs) break;
  }
  return false;
}

// Bounded wait; false (and *err set) when it gave up.  `bad` is a CTA flag in
// shared memory: once one wait of the CTA has given up, the later ones return
// at once (the ring is broken; the CTA finishes on invalid data, flagged).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err,
                                          volatile int* bad) {
  if (*bad) return false;
  if (mbar_poll(bar, parity)) return true;
  *bad = 1;
  if (err) atomicExch(err, kErrTimeout);
  return false;
}

// Bounded wait of a copy's own issuer for a copy that may still be in flight
// when the ring has broken: no error flag, no early return on `bad`; false when
// it gave up.
__device__ __forceinline__ bool mbar_drain(uint64_t* bar, uint32_t parity) {
  return mbar_poll(bar, parity);
}

// orders this thread's earlier generic-proxy accesses of shared memory
// before later async-proxy (TMA) writes to it
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 3-D tiled load of one box into shared memory, completing on `bar`
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace ns3d
