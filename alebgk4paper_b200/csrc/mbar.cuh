// mbar.cuh -- mbarrier and bulk-copy helpers shared by the sm_100a kernels
// (internal header).  Every wait is bounded: after kSpinLimit polls it gives
// up, marks the caller dead and returns, so a broken pipeline ends the kernel
// with an error bit instead of hanging the device.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace alebgk {

constexpr int kSpinLimit = 1 << 20;

__device__ __forceinline__ uint32_t smemAddr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbarInit(uint64_t *bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count));
}

// Makes barrier initialisation visible to the async proxy (TMA).
__device__ __forceinline__ void mbarInitFence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbarExpectTx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbarArrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(bar)) : "memory");
}

__device__ __forceinline__ bool mbarTryWait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smemAddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase.  A caller already marked dead does not
// wait again, so a broken pipeline costs one timeout, not one per stage.
__device__ __forceinline__ bool mbarWait(uint64_t *bar, uint32_t parity, bool &dead)
{
    if (dead) return false;
    for (int it = 0; it < kSpinLimit; ++it)
        if (mbarTryWait(bar, parity)) return true;
    dead = true;
    return false;
}

// Orders this thread's earlier generic-proxy accesses to shared memory before
// later async-proxy (bulk copy) accesses to it.
__device__ __forceinline__ void fenceProxyAsync()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One contiguous global -> shared copy through the bulk-copy engine; both
// addresses 16-byte aligned, bytes a multiple of 16.  Completes on bar.
__device__ __forceinline__ void bulkLoad(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1], %2, [%3];" ::"r"(smemAddr(dst)),
        "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smemAddr(bar))
        : "memory");
}

}  // namespace alebgk
