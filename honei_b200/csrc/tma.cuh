// Bulk (TMA) copies global -> shared with completion on an mbarrier, and a bounded
// wait for them.  No multicast: every copy lands in the issuing CTA's own shared
// memory.  The copy's addresses and size must be 16-byte aligned.
#pragma once

#include "hb2_common.cuh"

namespace hb2
{
    __device__ __forceinline__ uint32_t smem_addr(const void * p)
    {
        return (uint32_t)__cvta_generic_to_shared(p);
    }

    __device__ __forceinline__ void mbar_init(uint64_t * bar, unsigned count)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(bar)), "r"(count) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }

    __device__ __forceinline__ void mbar_expect_tx(uint64_t * bar, unsigned bytes)
    {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_addr(bar)), "r"(bytes)
                     : "memory");
    }

    __device__ __forceinline__ void bulk_g2s(void * dst, const void * src, unsigned bytes, uint64_t * bar)
    {
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
    }

    // init without the fences (several barriers initialised by one thread; the
    // caller fences once with mbar_init_fence)
    __device__ __forceinline__ void mbar_init_only(uint64_t * bar, unsigned count)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(bar)), "r"(count) : "memory");
    }

    __device__ __forceinline__ void mbar_init_fence()
    {
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }

    __device__ __forceinline__ bool mbar_try_wait(uint64_t * bar, unsigned parity)
    {
        uint32_t ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
        return ok != 0;
    }

    // bounded wait: false after limit_ns without completion
    __device__ __forceinline__ bool mbar_wait_bounded(uint64_t * bar, unsigned parity, unsigned long long limit_ns)
    {
        if (mbar_try_wait(bar, parity)) return true;
        unsigned long long t0 = global_ns();
        while (! mbar_try_wait(bar, parity))
            if (global_ns() - t0 > limit_ns) return false;
        return true;
    }
}
