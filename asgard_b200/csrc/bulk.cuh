// Shared-memory staging by the bulk-copy engine: mbarrier set-up, waits
// with a bound, and global -> shared copies (cp.async.bulk without
// multicast; the source is always this GPU's own memory).
#pragma once

#include <cstdint>

namespace asgk
{
namespace bulk
{
constexpr long long kWaitCycles = 1ll << 31; // about one second at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_init_fence()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar,
                                                      uint32_t bytes)
{
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

// a plain arrival: completes a phase that expects no copy
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(ok)
               : "r"(smem_u32(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}

// Waits until the phase with the given parity has completed, or gives up
// after kWaitCycles.  The decision is warp-uniform.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar,
                                                  uint32_t parity)
{
  long long const t0 = clock64();
  while (true)
  {
    bool const ok = mbar_try_wait(bar, parity);
    if (__all_sync(0xffffffffu, ok))
      return true;
    if (__any_sync(0xffffffffu, clock64() - t0 > kWaitCycles))
      return false;
  }
}

// global -> shared bulk copy (no multicast), completion counted on bar;
// both addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src,
                                         uint32_t bytes, uint64_t *bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::"
               "bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// orders this thread's earlier shared-memory accesses before later
// async-proxy (bulk copy) accesses
__device__ __forceinline__ void fence_proxy_async_smem()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
} // namespace bulk
} // namespace asgk
