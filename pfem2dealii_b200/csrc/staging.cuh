// Bulk asynchronous copies global -> shared memory (cp.async.bulk, the TMA
// engine's 1D form) completed through an mbarrier, with bounded waits.
//
// Rules kept here: source and destination 16-byte aligned, sizes multiples of
// 16 bytes, no multicast; every wait gives up after a fixed number of polls
// and reports it, so a kernel can never hang on a copy.
#pragma once

#include <cstdint>

namespace pfem2 {

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make initialised barriers visible to the async proxy.
__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Order this thread's earlier shared-memory accesses (generic proxy) before
// later bulk copies into the same buffer (async proxy).
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

constexpr uint32_t MBAR_POLL_LIMIT = 1u << 22;

// Wait for phase `parity` of the barrier; false after MBAR_POLL_LIMIT polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    for (uint32_t k = 0; k < MBAR_POLL_LIMIT; ++k) {
        if (mbar_test(bar, parity)) return true;
        if (k > 16) __nanosleep(32);
    }
    return false;
}

}  // namespace pfem2
