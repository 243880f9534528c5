// s2d_async.cuh -- TMA bulk copies (cp.async.bulk) into shared memory with mbarrier
// completion, and a bounded wait.
//
// Used to stage whole contiguous rows (state rows, forcing rows) into shared
// memory at kernel start so that their HBM/L2 latency overlaps the row FFT
// that precedes their use.  No cluster multicast anywhere.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace s2d {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// make the initialised barrier visible to the async (TMA) proxy
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// bytes (multiple of 16, both addresses 16-byte aligned) global -> this CTA's shared memory
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// nanoseconds of the GPU's global timer
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// default limit of a device-side wait: far above any legitimate wait in these kernels
// (a bulk copy or an MMA group of microseconds), short enough that a wait that can never
// end returns well inside a host-side timeout
constexpr uint64_t kWaitLimitNs = 50ull * 1000ull * 1000ull;   // 50 ms

// Wait for phase `parity` of the barrier for at most `limit_ns` of global-timer time.
// On giving up, records `code` in the device error word and returns false; the
// caller's results are then invalid and the host reports the error at its next
// synchronization (s2d_synchronize / any call that reads the error word).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err, int code,
                                                  uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (globaltimer_ns() - t0 > limit_ns) break;
  }
  if (err) atomicExch(err, code);
  return false;
}

}  // namespace s2d
