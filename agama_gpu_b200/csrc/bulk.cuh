// bulk.cuh -- bulk (TMA) copies from global to shared memory with an mbarrier.
//
// One thread of the block arms the barrier with the byte count and issues
// cp.async.bulk; every thread then waits for the barrier's phase.  The copy is
// untiled: source and destination 16-byte aligned, size a multiple of 16 bytes
// (callers copy whole 32-byte FP32 records).  Waits are bounded: a wait that
// gives up returns false and the caller falls back to reading global memory.
#pragma once
#include <stdint.h>

__device__ __forceinline__ unsigned smem_addr(const void* p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(bar)), "r"(count)
                 : "memory");
    // make the initialised barrier visible to the async proxy (the bulk copies)
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// before an async-proxy write to shared memory that generic loads read earlier
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// one arrival that also expects `bytes` of transactions on the barrier
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes,
                                              uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                 "[%0], [%1], %2, [%3];"
                 :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// wait for the barrier's phase `parity` to complete, at most `tries` polls
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, int tries)
{
    for (int i = 0; i < tries; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
