// Bulk asynchronous copies (the TMA engine) and shared-memory mbarriers for
// the pipelined Born kernels, in inline PTX for sm_100a.
//
// Only plain global -> shared bulk copies are used (no cluster multicast):
// the copies read this GPU's own memory.  Every wait is bounded: after
// ~2^31 clock cycles (about a second at the B200's clocks) without the
// barrier completing, the waiting thread reports a timeout and the kernel
// abandons its work (the host reads the fault word and fails the call).
#pragma once

#include <stdint.h>

#include <atomic>

namespace odt {

// Default bound of every mbarrier wait: 2^31 clock cycles (about a second).
// The steady waits of the pipelined Born kernels take the handle's limit
// instead (ODT_WAIT_LIMIT_CYCLES at odt_create); the waits that drain a
// CTA's copies in flight before it gives up always keep this one, so no bulk
// copy is still writing shared memory when the CTA exits.
constexpr long long kWaitLimitCycles = 1LL << 31;

#if defined(__CUDA_ARCH__)

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// make barrier initialisation visible to the async proxy (the copy engine)
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// order this thread's earlier generic-proxy accesses of shared memory before
// later async-proxy accesses (a bulk copy about to overwrite a buffer)
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// global -> shared bulk copy of `bytes` (multiple of 16, both addresses
// 16-byte aligned), completing `bytes` transactions on `bar`
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// One non-blocking poll of phase `parity` of `bar`.
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for phase `parity` of `bar`; false once `limit` clock cycles
// have passed without the phase completing.  A limit of 0 is one
// non-blocking poll (try_wait itself may suspend the thread for a while).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit = kWaitLimitCycles) {
  if (limit <= 0) return mbar_test_wait(bar, parity);
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return false;
  }
  return true;
}

// *p += v component-wise in L2 (red.global.add.v2.f32: round to nearest;
// subnormal inputs and results flush to zero, which the Born fields never
// reach), with no value returned, so the thread does not wait for it: the
// steady Born passes accumulate Field this way
__device__ __forceinline__ void red_add2(float2* p, float2 v) {
  asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(v.x), "f"(v.y) : "memory");
}

#endif  // __CUDA_ARCH__

// Host side: one flag per (kernel instantiation, device) saying that the
// kernel's dynamic shared-memory limit has been raised on that device.
struct DeviceFlags {
  std::atomic<unsigned long long> bits{0};
  bool test(int dev) const { return dev < 64 && ((bits.load() >> dev) & 1ull); }
  void set(int dev) {
    if (dev < 64) bits.fetch_or(1ull << dev);
  }
};

// fault codes written by the pipelined kernels (first one wins)
enum PipeFault { kFaultNone = 0, kFaultTimeout = 1, kFaultAlign = 2 };

}  // namespace odt
