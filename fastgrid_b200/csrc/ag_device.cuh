// Shared device-side helpers: PTX wrappers for the TMA bulk-copy engine and
// mbarriers, bounded waits, and the error-status word kernels report through.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace agd {

// Error bits a kernel may set in its status word (read back by the host).
enum : unsigned {
  ST_WAIT_TIMEOUT = 1u,   // a bounded mbarrier wait gave up
  ST_BAD_INPUT = 2u,      // an index or size outside the launch's stated bounds
};

constexpr long long kWaitLimit = 1ll << 26;  // polls before a wait gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Arrive on `bar` and announce `bytes` of incoming asynchronous transfer.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// One 1-D bulk copy global -> shared, completion signalled on `bar`.
// dst, src 16-byte aligned; bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for phase `parity` of `bar` to complete, at most kWaitLimit polls.
// Returns false (and sets ST_WAIT_TIMEOUT in *status) if it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, unsigned* status) {
  for (long long i = 0; i < kWaitLimit; i++)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(status, ST_WAIT_TIMEOUT);
  return false;
}

// The same with an explicit poll limit (a test hook uses a few polls on a
// barrier nothing arrives on, to make the expiry path run).
__device__ __forceinline__ bool mbar_wait_limit(uint64_t* bar, unsigned parity, unsigned* status, int limit) {
  for (int i = 0; i < limit; i++)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(status, ST_WAIT_TIMEOUT);
  return false;
}

__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

}  // namespace agd
