// bulk.cuh -- bulk-async (TMA engine) copies into shared memory, completed on
// an mbarrier, and the bounded wait used on them.
//
// cp.async.bulk moves a contiguous global range into this CTA's shared memory
// without a register round trip; the copy engine signals its bytes on an
// mbarrier whose phase completes when the expected byte count has arrived.
// Every wait here has a time limit: a phase that does not complete (a byte
// count declared but never delivered) makes the wait return false instead of
// spinning forever, and the kernel reports that through a status word.
// Loads are plain (no cluster multicast): the source is this GPU's memory.
#pragma once
#include <stdint.h>

namespace zk {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Makes initialised barriers visible to the copy engine (async proxy).
__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Orders this thread's earlier generic-proxy accesses of shared memory before
// later bulk copies into it.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// One arrival that also raises the phase's expected byte count by tx.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t tx)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(tx) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of the given parity to complete, for at most limit_ns
// of GPU time; false if it did not.  The barrier is tested once more after the
// limit, so a CTA that was descheduled past it does not report a false timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint64_t limit_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > limit_ns) return mbar_try_wait(bar, parity);
    }
}

// bytes from global src to shared dst, signalled on bar; dst, src and bytes
// are multiples of 16.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

}  // namespace zk
